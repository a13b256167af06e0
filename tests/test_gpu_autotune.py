"""Launch shapes and the autotuner (eimp_b200/autotune.py): every launch shape
of the dosage kernel, the match search and the persistent beam gives the same
outputs bit for bit, the tuner leaves one of the candidates set, and invalid
shapes are refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_launch_shapes_do_not_change_results():
    import torch
    from eimp_b200 import synth
    from eimp_b200._lib import EimpError
    from eimp_b200.autotune import KNOBS, get, set_shape, tune_group
    from eimp_b200.batch import DensityGroup
    from eimp_b200.engine import PhaseParams
    panel, groups = synth.generate("cfg1")
    tg = groups[0]
    dev = torch.device("cuda", 0)
    d_full = torch.from_numpy(panel.sitemajor.view(np.int64)).to(dev)
    d_af = torch.from_numpy(panel.af.astype(np.float32)).to(dev)
    hm, sm, cm = synth.typed_views(panel, tg.typed)
    g = DensityGroup(0, d_full, d_af, panel.nhaps, tg.typed, hm, sm, cm, tg.gt[:40], PhaseParams(K=1024, beamwidth=64),
                     batch_targets=16)
    g.enqueue()
    g.ctx.synchronize()
    ref = [x.clone() for x in (g.d_mats, g.d_pats, g.d_pdm, g.d_dos, g.d_bits)]
    for k, (_, vals) in KNOBS.items():
        for v in vals:
            set_shape(g, k, v)
            assert get(g, k) == v
            for x in (g.d_mats, g.d_dos, g.d_bits):
                x.zero_()
            g.enqueue()
            g.ctx.synchronize()
            for a, b in zip((g.d_mats, g.d_pats, g.d_pdm, g.d_dos, g.d_bits), ref):
                assert torch.equal(a, b), (k, v)
        set_shape(g, k, vals[0])
    with pytest.raises(EimpError):
        set_shape(g, "dosage_span", 5)
    res = tune_group(g, reps=1)
    for k, r in res.items():
        assert r["chosen"] in KNOBS[k][1] and get(g, k) == r["chosen"]
    for a, b in zip((g.d_mats, g.d_pats, g.d_pdm, g.d_dos, g.d_bits), ref):
        assert torch.equal(a, b)
    g.close()
