"""GPU parity: phasing with start phases carried over from a previous chunk
(VCFData::getStartPhase, Target.cpp:311-312, 443) against the reference's own
Target::phase (oracle/_ref) with the same chunkStartPhase, with and without
pre-phasing; bit-exact."""
import numpy as np
import pytest

from conftest import golden_path

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prephase", [False, True])
def test_start_phases_vs_reference(ctx, prephase):
    from eimp_b200.engine import PhaseParams, Phaser
    from oracle import refcore
    if not refcore.available():
        pytest.skip("reference sources not compiled (oracle/_ref)")
    g = np.load(golden_path("golden_tiny.npz"))
    hm, sm, cm, gt = g["hapmajor_typed"], g["sitemajor_typed"], g["cm_typed"], g["gt"]
    n = gt.shape[0]
    phases = (np.arange(n) % 3 != 0).astype(np.uint8)   # mixed Ref / Alt starts
    ph = Phaser(ctx, hm, sm, cm)
    ph.setStartPhases(phases)
    got = ph.phase(PhaseParams(K=64, beamwidth=16, doPrePhasing=prephase), gt)
    base = None
    ph.setStartPhases(None)
    base = ph.phase(PhaseParams(K=64, beamwidth=16, doPrePhasing=prephase), gt)
    rc = refcore.RefCore.typed_only(hm, sm, cm, gt, g["af_full"][g["typed"]])
    rc.set_start_phases(phases)
    rc.set_params(refcore.PhaseParams(K=64, beamwidth=16, doPrePhasing=prephase))
    ref = [rc.phase(t) for t in range(n)]
    rc.close()
    for t in range(n):
        for name, a, b in zip(("mat", "pat", "dm", "dp"), [x[t] for x in got[:4]], ref[t][:4]):
            np.testing.assert_array_equal(a, b, err_msg=f"target {t} {name}")
        assert got[4][t] == np.float32(ref[t][4]) and got[5][t] == ref[t][5]
    # an Alt start changes the phased haplotypes of the targets it is given to
    assert any(not np.array_equal(got[0][t], base[0][t]) for t in range(n) if phases[t])
