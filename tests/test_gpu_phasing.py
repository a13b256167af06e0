"""GPU parity: beam phasing (Target::phase) against the golden fixtures made by
the reference and against the oracle restatement.  Phased haplotypes must be
bit-exact; phasing dosages and confidences are floats computed in the
reference's operation order and are compared exactly as well (tolerance 0)."""
import numpy as np
import pytest

from conftest import golden_path
from eimp_b200.bits import W, unpack_rows

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    return np.load(golden_path("golden_tiny.npz"))


def first_diff(a, b, M):
    ua, ub = unpack_rows(a, M), unpack_rows(b, M)
    d = np.nonzero(ua != ub)[0]
    return d[:5]


@pytest.mark.parametrize("K", [64, 50, 200])
def test_phase_golden(ctx, g, K):
    from eimp_b200.engine import PhaseParams, Phaser
    pre = f"K{K}_"
    ph = Phaser(ctx, g["hapmajor_typed"], g["sitemajor_typed"], g["cm_typed"])
    mats, pats, dm, dp, tc, nc = ph.phase(PhaseParams(K=K, beamwidth=16), g["gt"])
    M = int(g["M"])
    for t in range(g["gt"].shape[0]):
        assert np.array_equal(mats[t], g[pre + "mat"][t]), (t, first_diff(mats[t], g[pre + "mat"][t], M))
        assert np.array_equal(pats[t], g[pre + "pat"][t]), t
        np.testing.assert_array_equal(dm[t], g[pre + "dos_mat"][t])
        np.testing.assert_array_equal(dp[t], g[pre + "dos_pat"][t])
    np.testing.assert_array_equal(tc, g[pre + "totalconf"])
    np.testing.assert_array_equal(nc, g[pre + "ncallsites"])


@pytest.mark.parametrize("prephase,beam", [(False, 32), (True, 32), (True, 4)])
def test_phase_vs_oracle_smalltest(ctx, smalltest, prephase, beam):
    """beam 4: most prunes keep the 4 best of more candidates."""
    from eimp_b200.engine import PhaseParams, Phaser
    from eimp_b200.synth import typed_views
    from oracle import restate as R
    panel, groups = smalltest
    tg = groups[0]
    hm, sm, cm = typed_views(panel, tg.typed)
    ph = Phaser(ctx, hm, sm, cm)
    pp = PhaseParams(K=200, beamwidth=beam, doPrePhasing=prephase)
    mats, pats, dm, dp, tc, nc = ph.phase(pp, tg.gt)
    P = R.params_c(K=200, beamwidth=beam, doPrePhasing=prephase)
    om, op, odm, odp = R.phase_many(tg.gt, hm, sm, cm, P, 8)
    for t in range(tg.gt.shape[0]):
        assert np.array_equal(mats[t], om[t]), (t, first_diff(mats[t], om[t], len(tg.typed)))
        assert np.array_equal(pats[t], op[t]), t
        np.testing.assert_array_equal(dm[t], odm[t])
        np.testing.assert_array_equal(dp[t], odp[t])


def test_phase_vs_oracle_cfg1_sample(ctx):
    """cfg1 (5000 haplotypes, 2000 typed sites, K=1024, beam 64): 24 targets."""
    from eimp_b200 import synth
    from eimp_b200.engine import PhaseParams, Phaser
    from eimp_b200.synth import typed_views
    from oracle import restate as R
    panel, groups = synth.generate("cfg1")
    tg = groups[0]
    nt = 24
    hm, sm, cm = typed_views(panel, tg.typed)
    ph = Phaser(ctx, hm, sm, cm)
    mats, pats, dm, dp, tc, nc = ph.phase(PhaseParams(K=1024, beamwidth=64), tg.gt[:nt])
    om, op, odm, odp = R.phase_many(tg.gt[:nt], hm, sm, cm, R.params_c(K=1024, beamwidth=64), 8)
    bad = [t for t in range(nt) if not (np.array_equal(mats[t], om[t]) and np.array_equal(pats[t], op[t])
                                        and np.array_equal(dm[t], odm[t]) and np.array_equal(dp[t], odp[t]))]
    assert not bad, f"targets differing from the oracle: {bad}"
